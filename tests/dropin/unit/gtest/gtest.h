// gtest/gtest.h -- the subset of GoogleTest's test macros that the
// reference's unit tests of this path use (TEST, EXPECT_/ASSERT_ EQ NE LT LE
// GT GE NEAR TRUE FALSE THROW, EXPECT_DOUBLE_EQ / FLOAT_EQ, GTEST_SKIP,
// streamed messages), so those test files
// compile unchanged here without GoogleTest.  Test infrastructure only.
//
// Each TEST registers a function; tests/dropin/unit/gtest_main.cpp runs
// them in order (optionally filtered), prints one "[ RUN ]" line and one of
// "[ OK ]", "[ FAILED ]", "[ SKIPPED ]" per test, and exits non-zero if any
// failed.  An exception escaping a test fails it.
#pragma once

#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <functional>
#include <sstream>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace gtest_shim {

struct TestCase {
  std::string suite, name;
  void (*fn)();
};

inline std::vector<TestCase>& registry() {
  static std::vector<TestCase> r;
  return r;
}

struct State {
  bool failed = false;
  bool skipped = false;
};
inline State& state() {
  static State s;
  return s;
}

struct Registrar {
  Registrar(const char* suite, const char* name, void (*fn)()) {
    registry().push_back(TestCase{suite, name, fn});
  }
};

class Message {
 public:
  template <class T>
  Message& operator<<(const T& v) {
    s_ << v;
    return *this;
  }
  std::string str() const { return s_.str(); }

 private:
  std::ostringstream s_;
};

// `helper = Message() << ...;` reports when the assignment runs (after the
// streamed message is complete); returns void so `return helper = ...;`
// leaves a test body after a fatal failure.
struct FailureHelper {
  const char* file;
  int line;
  std::string what;
  void operator=(const Message& m) const {
    state().failed = true;
    std::printf("%s:%d: Failure\n%s\n%s\n", file, line, what.c_str(), m.str().c_str());
  }
};

struct SkipHelper {
  void operator=(const Message& m) const {
    state().skipped = true;
    const std::string s = m.str();
    if (!s.empty()) std::printf("Skipped: %s\n", s.c_str());
  }
};

struct Result {
  bool ok;
  std::string what;
  explicit operator bool() const { return ok; }
};

template <class T, class = void>
struct Streamable : std::false_type {};
template <class T>
struct Streamable<T, std::void_t<decltype(std::declval<std::ostream&>() << std::declval<const T&>())>>
    : std::true_type {};

template <class T, class = void>
struct HasSize : std::false_type {};
template <class T>
struct HasSize<T, std::void_t<decltype(std::declval<const T&>().size())>> : std::true_type {};

// The value in a failure message; enums print their integer, containers
// their size, other values without an output operator a placeholder.
template <class T>
std::string show(const T& v) {
  std::ostringstream s;
  s.precision(17);
  if constexpr (std::is_enum_v<T>)
    s << static_cast<long long>(v);
  else if constexpr (Streamable<T>::value)
    s << v;
  else if constexpr (HasSize<T>::value)
    s << "{container of " << v.size() << " elements}";
  else
    s << "{value}";
  return s.str();
}

template <class A, class B, class Op>
Result compare(const A& a, const B& b, Op op, const char* macro, const char* ea, const char* eb) {
  if (op(a, b)) return Result{true, {}};
  return Result{false, std::string(macro) + "(" + ea + ", " + eb + ")\n  left:  " + show(a) +
                           "\n  right: " + show(b)};
}

template <class A, class B, class C>
Result near(const A& a, const B& b, const C& tol, const char* ea, const char* eb, const char* et) {
  const double d = std::fabs(static_cast<double>(a) - static_cast<double>(b));
  if (d <= static_cast<double>(tol)) return Result{true, {}};
  return Result{false, std::string("EXPECT_NEAR(") + ea + ", " + eb + ", " + et +
                           ")\n  difference " + show(d) + " exceeds " +
                           show(static_cast<double>(tol)) + "\n  left:  " + show(a) +
                           "\n  right: " + show(b)};
}

// Within 4 units in the last place, GoogleTest's floating-point equality.
template <class T>
Result ulp_eq(T a, T b, const char* macro, const char* ea, const char* eb) {
  static_assert(std::is_floating_point_v<T>);
  using U = std::conditional_t<sizeof(T) == 8, long long, int>;
  auto key = [](T x) {
    U u;
    std::memcpy(&u, &x, sizeof u);
    return u < 0 ? std::numeric_limits<U>::min() - u : u;  // sign-magnitude -> ordered
  };
  bool ok = a == b;
  if (!ok && !std::isnan(a) && !std::isnan(b)) {
    const U ka = key(a), kb = key(b);
    ok = (ka > kb ? ka - kb : kb - ka) <= 4;
  }
  if (ok) return Result{true, {}};
  return Result{false, std::string(macro) + "(" + ea + ", " + eb + ")\n  left:  " + show(a) +
                           "\n  right: " + show(b)};
}

inline Result truth(bool v, bool want, const char* macro, const char* e) {
  if (v == want) return Result{true, {}};
  return Result{false, std::string(macro) + "(" + e + ")"};
}

}  // namespace gtest_shim

#define TDMD_GT_CONCAT2_(a, b) a##b
#define TDMD_GT_CONCAT_(a, b) TDMD_GT_CONCAT2_(a, b)
#define TDMD_GT_NAME_(suite, name) TDMD_GT_CONCAT_(gtest_case_##suite##_, name)

#define TEST(suite, name)                                                               \
  static void TDMD_GT_NAME_(suite, name)();                                             \
  static ::gtest_shim::Registrar TDMD_GT_CONCAT_(TDMD_GT_NAME_(suite, name), _reg_)(    \
      #suite, #name, &TDMD_GT_NAME_(suite, name));                                      \
  static void TDMD_GT_NAME_(suite, name)()

#define TDMD_GT_FAIL_(what) ::gtest_shim::FailureHelper{__FILE__, __LINE__, (what)} = ::gtest_shim::Message()

#define TDMD_GT_EXPECT_(result) \
  if (const ::gtest_shim::Result tdmd_gt_r_ = (result)) {                               \
  } else                                                                                \
    TDMD_GT_FAIL_(tdmd_gt_r_.what)

#define TDMD_GT_ASSERT_(result) \
  if (const ::gtest_shim::Result tdmd_gt_r_ = (result)) {                               \
  } else                                                                                \
    return TDMD_GT_FAIL_(tdmd_gt_r_.what)

#define TDMD_GT_CMP_(a, b, op, macro) \
  ::gtest_shim::compare((a), (b), [](const auto& x, const auto& y) { return x op y; }, macro, #a, #b)

#define EXPECT_EQ(a, b) TDMD_GT_EXPECT_(TDMD_GT_CMP_(a, b, ==, "EXPECT_EQ"))
#define EXPECT_NE(a, b) TDMD_GT_EXPECT_(TDMD_GT_CMP_(a, b, !=, "EXPECT_NE"))
#define EXPECT_LT(a, b) TDMD_GT_EXPECT_(TDMD_GT_CMP_(a, b, <, "EXPECT_LT"))
#define EXPECT_LE(a, b) TDMD_GT_EXPECT_(TDMD_GT_CMP_(a, b, <=, "EXPECT_LE"))
#define EXPECT_GT(a, b) TDMD_GT_EXPECT_(TDMD_GT_CMP_(a, b, >, "EXPECT_GT"))
#define EXPECT_GE(a, b) TDMD_GT_EXPECT_(TDMD_GT_CMP_(a, b, >=, "EXPECT_GE"))
#define ASSERT_EQ(a, b) TDMD_GT_ASSERT_(TDMD_GT_CMP_(a, b, ==, "ASSERT_EQ"))
#define ASSERT_NE(a, b) TDMD_GT_ASSERT_(TDMD_GT_CMP_(a, b, !=, "ASSERT_NE"))
#define ASSERT_LT(a, b) TDMD_GT_ASSERT_(TDMD_GT_CMP_(a, b, <, "ASSERT_LT"))
#define ASSERT_LE(a, b) TDMD_GT_ASSERT_(TDMD_GT_CMP_(a, b, <=, "ASSERT_LE"))
#define ASSERT_GT(a, b) TDMD_GT_ASSERT_(TDMD_GT_CMP_(a, b, >, "ASSERT_GT"))
#define ASSERT_GE(a, b) TDMD_GT_ASSERT_(TDMD_GT_CMP_(a, b, >=, "ASSERT_GE"))
#define EXPECT_NEAR(a, b, tol) TDMD_GT_EXPECT_(::gtest_shim::near((a), (b), (tol), #a, #b, #tol))
#define ASSERT_NEAR(a, b, tol) TDMD_GT_ASSERT_(::gtest_shim::near((a), (b), (tol), #a, #b, #tol))
#define EXPECT_TRUE(c) TDMD_GT_EXPECT_(::gtest_shim::truth(static_cast<bool>(c), true, "EXPECT_TRUE", #c))
#define EXPECT_FALSE(c) TDMD_GT_EXPECT_(::gtest_shim::truth(static_cast<bool>(c), false, "EXPECT_FALSE", #c))
#define ASSERT_TRUE(c) TDMD_GT_ASSERT_(::gtest_shim::truth(static_cast<bool>(c), true, "ASSERT_TRUE", #c))
#define ASSERT_FALSE(c) TDMD_GT_ASSERT_(::gtest_shim::truth(static_cast<bool>(c), false, "ASSERT_FALSE", #c))
#define EXPECT_DOUBLE_EQ(a, b) \
  TDMD_GT_EXPECT_(::gtest_shim::ulp_eq<double>((a), (b), "EXPECT_DOUBLE_EQ", #a, #b))
#define EXPECT_FLOAT_EQ(a, b) \
  TDMD_GT_EXPECT_(::gtest_shim::ulp_eq<float>((a), (b), "EXPECT_FLOAT_EQ", #a, #b))
#define TDMD_GT_THROWS_(stmt, type, fatal_return)                                      \
  if (const ::gtest_shim::Result tdmd_gt_r_ = [&] {                                    \
        try {                                                                          \
          stmt;                                                                        \
        } catch (const type&) {                                                        \
          return ::gtest_shim::Result{true, {}};                                       \
        } catch (...) {                                                                \
          return ::gtest_shim::Result{false, "EXPECT_THROW(" #stmt ", " #type           \
                                             "): threw another type"};                 \
        }                                                                              \
        return ::gtest_shim::Result{false, "EXPECT_THROW(" #stmt ", " #type            \
                                           "): did not throw"};                        \
      }()) {                                                                           \
  } else                                                                               \
    fatal_return TDMD_GT_FAIL_(tdmd_gt_r_.what)
#define EXPECT_THROW(stmt, type) TDMD_GT_THROWS_(stmt, type, )
#define ASSERT_THROW(stmt, type) TDMD_GT_THROWS_(stmt, type, return)
#define GTEST_SKIP() return ::gtest_shim::SkipHelper{} = ::gtest_shim::Message()
#define FAIL() return TDMD_GT_FAIL_("FAIL()")
#define ADD_FAILURE() TDMD_GT_FAIL_("ADD_FAILURE()")
