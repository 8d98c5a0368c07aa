// A minimal stand-in for <gtest/gtest.h> (GoogleTest is not installed here),
// enough to compile and run the reference's scheduler tests unchanged:
// TEST, TEST_F, ::testing::Test with SetUp/TearDown, the ASSERT_/EXPECT_
// comparison macros with `<< message` streaming, and GTEST_SKIP().
// ASSERT_* failures end the test (an exception caught by the runner);
// EXPECT_* failures are recorded and the test continues.  run_all() runs
// every registered test and returns 0 only if none failed.
//
// This is test infrastructure: it lets the reference's own tests check the
// B200 engine's schedule_pairhmm through the unchanged symbol.
#pragma once
#include <cmath>
#include <cstdio>
#include <functional>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

namespace testing {
class Test {
 public:
  virtual ~Test() = default;
  virtual void SetUp() {}
  virtual void TearDown() {}
  virtual void TestBody() = 0;
};
}  // namespace testing

namespace gtm {

struct FatalFailure {};
struct Skipped {};

struct Registry {
  struct Entry {
    std::string name;
    std::function<testing::Test*()> make;
  };
  std::vector<Entry> tests;
  std::vector<std::string> traces;  // SCOPED_TRACE messages in scope
  int failures_in_test = 0;
  static Registry& get() {
    static Registry r;
    return r;
  }
};

inline int add_test(const char* suite, const char* name, std::function<testing::Test*()> make) {
  Registry::get().tests.push_back({std::string(suite) + "." + name, std::move(make)});
  return 0;
}

template <class T>
std::string show(const T& v) {
  if constexpr (std::is_arithmetic<T>::value || std::is_same<T, std::string>::value) {
    std::ostringstream s;
    s.precision(17);
    s << v;
    return s.str();
  } else {
    return "<value>";
  }
}

// Reports a failure when it goes out of scope, with any streamed message;
// a fatal one then throws to end the test.
class Failure {
 public:
  Failure(bool fatal, const char* file, int line, std::string what)
      : fatal_(fatal), file_(file), line_(line), what_(std::move(what)) {}
  template <class T>
  Failure& operator<<(const T& v) {
    msg_ << v;
    return *this;
  }
  ~Failure() noexcept(false) {
    std::fprintf(stderr, "%s:%d: Failure\n%s\n%s\n", file_, line_, what_.c_str(),
                 msg_.str().c_str());
    for (const std::string& t : Registry::get().traces) std::fprintf(stderr, "  trace: %s\n", t.c_str());
    Registry::get().failures_in_test++;
    if (fatal_) throw FatalFailure{};
  }

 private:
  bool fatal_;
  const char* file_;
  int line_;
  std::string what_;
  std::ostringstream msg_;
};

class Skip {
 public:
  Skip(const char* file, int line) : file_(file), line_(line) {}
  template <class T>
  Skip& operator<<(const T& v) {
    msg_ << v;
    return *this;
  }
  ~Skip() noexcept(false) {
    std::fprintf(stderr, "%s:%d: Skipped\n%s\n", file_, line_, msg_.str().c_str());
    throw Skipped{};
  }

 private:
  const char* file_;
  int line_;
  std::ostringstream msg_;
};

class ScopedTrace {
 public:
  template <class T>
  ScopedTrace(const char* file, int line, const T& msg) {
    std::ostringstream s;
    s << file << ":" << line << ": " << msg;
    Registry::get().traces.push_back(s.str());
  }
  ~ScopedTrace() { Registry::get().traces.pop_back(); }
};

template <class A, class B>
std::string cmp_text(const char* op, const char* ea, const char* eb, const A& a, const B& b) {
  return std::string("Expected: (") + ea + ") " + op + " (" + eb + "), actual: " + show(a) +
         " vs " + show(b);
}

inline int run_all() {
  Registry& r = Registry::get();
  int failed = 0, skipped = 0, passed = 0;
  for (auto& t : r.tests) {
    std::printf("[ RUN      ] %s\n", t.name.c_str());
    std::fflush(stdout);
    r.failures_in_test = 0;
    r.traces.clear();
    bool skip = false;
    testing::Test* obj = t.make();
    try {
      obj->SetUp();
      obj->TestBody();
    } catch (const FatalFailure&) {
    } catch (const Skipped&) {
      skip = true;
    } catch (const std::exception& e) {
      std::fprintf(stderr, "uncaught exception: %s\n", e.what());
      r.failures_in_test++;
    }
    try {
      obj->TearDown();
    } catch (...) {
      r.failures_in_test++;
    }
    delete obj;
    if (r.failures_in_test) {
      ++failed;
      std::printf("[  FAILED  ] %s\n", t.name.c_str());
    } else if (skip) {
      ++skipped;
      std::printf("[  SKIPPED ] %s\n", t.name.c_str());
    } else {
      ++passed;
      std::printf("[       OK ] %s\n", t.name.c_str());
    }
    std::fflush(stdout);
  }
  std::printf("[==========] %zu tests: %d passed, %d skipped, %d failed\n", r.tests.size(), passed,
              skipped, failed);
  return failed ? 1 : 0;
}

}  // namespace gtm

#define GTM_CLASS(suite, name) suite##_##name##_Test
#define GTM_DEFINE(suite, name, base)                                                     \
  class GTM_CLASS(suite, name) : public base {                                            \
   public:                                                                                \
    void TestBody() override;                                                             \
  };                                                                                      \
  static int gtm_reg_##suite##_##name = ::gtm::add_test(                                  \
      #suite, #name, [] { return static_cast<::testing::Test*>(new GTM_CLASS(suite, name)); }); \
  void GTM_CLASS(suite, name)::TestBody()
#define TEST(suite, name) GTM_DEFINE(suite, name, ::testing::Test)
#define TEST_F(fixture, name) GTM_DEFINE(fixture, name, fixture)

#define GTM_CHECK(cond, fatal, text) \
  if (cond)                          \
    ;                                \
  else                               \
    ::gtm::Failure(fatal, __FILE__, __LINE__, text)

#define GTM_CMP(a, b, op, fatal) \
  GTM_CHECK((a)op(b), fatal, ::gtm::cmp_text(#op, #a, #b, (a), (b)))

#define ASSERT_TRUE(c) GTM_CHECK(static_cast<bool>(c), true, "Expected true: " #c)
#define ASSERT_FALSE(c) GTM_CHECK(!static_cast<bool>(c), true, "Expected false: " #c)
#define EXPECT_TRUE(c) GTM_CHECK(static_cast<bool>(c), false, "Expected true: " #c)
#define EXPECT_FALSE(c) GTM_CHECK(!static_cast<bool>(c), false, "Expected false: " #c)
#define ASSERT_EQ(a, b) GTM_CMP(a, b, ==, true)
#define ASSERT_NE(a, b) GTM_CMP(a, b, !=, true)
#define ASSERT_LT(a, b) GTM_CMP(a, b, <, true)
#define ASSERT_LE(a, b) GTM_CMP(a, b, <=, true)
#define ASSERT_GT(a, b) GTM_CMP(a, b, >, true)
#define ASSERT_GE(a, b) GTM_CMP(a, b, >=, true)
#define EXPECT_EQ(a, b) GTM_CMP(a, b, ==, false)
#define EXPECT_NE(a, b) GTM_CMP(a, b, !=, false)
#define EXPECT_LT(a, b) GTM_CMP(a, b, <, false)
#define EXPECT_LE(a, b) GTM_CMP(a, b, <=, false)
#define EXPECT_GT(a, b) GTM_CMP(a, b, >, false)
#define EXPECT_GE(a, b) GTM_CMP(a, b, >=, false)
#define GTM_NEAR(a, b, tol, fatal)                                                        \
  GTM_CHECK(std::fabs(static_cast<double>(a) - static_cast<double>(b)) <=                 \
                static_cast<double>(tol),                                                 \
            fatal,                                                                        \
            std::string("Expected |" #a " - " #b "| <= " #tol ", actual: ") +             \
                ::gtm::show(static_cast<double>(a)) + " vs " +                            \
                ::gtm::show(static_cast<double>(b)))
#define ASSERT_NEAR(a, b, tol) GTM_NEAR(a, b, tol, true)
#define EXPECT_NEAR(a, b, tol) GTM_NEAR(a, b, tol, false)
#define GTEST_SKIP() ::gtm::Skip(__FILE__, __LINE__)
#define GTM_CAT2(a, b) a##b
#define GTM_CAT(a, b) GTM_CAT2(a, b)
#define SCOPED_TRACE(msg) ::gtm::ScopedTrace GTM_CAT(gtm_trace_, __LINE__)(__FILE__, __LINE__, (msg))
