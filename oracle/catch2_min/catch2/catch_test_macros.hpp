// catch_test_macros.hpp - a minimal test runner exposing the Catch2 v3 macro
// names that the reference project's test files use (TEST_CASE, CHECK, REQUIRE,
// CHECK_FALSE, REQUIRE_FALSE, CHECK_THROWS_AS, REQUIRE_THROWS_AS, CHECK_NOTHROW,
// INFO, SKIP, SUCCEED, FAIL), so that those files compile unchanged without the
// Catch2 library (which the reference fetches over the network at configure
// time). Test infrastructure: it links with catch_main.cpp.
//
// Semantics kept from Catch2: CHECK records a failure and continues, REQUIRE
// records it and ends the test case, SKIP ends the test case as skipped, a
// stray exception fails the test case. Expressions are reported as written (no
// operand decomposition).
#pragma once

#include <cstdio>
#include <exception>
#include <sstream>
#include <string>
#include <vector>

namespace catch_min {

struct TestCase {
  const char* name;
  const char* tags;
  void (*fn)();
};

inline std::vector<TestCase>& registry() {
  static std::vector<TestCase> r;
  return r;
}

struct Registrar {
  Registrar(const char* name, const char* tags, void (*fn)()) { registry().push_back({name, tags, fn}); }
};

struct State {
  int failures = 0;      // failed assertions in the current test case
  long assertions = 0;   // all assertions in the run
  std::vector<std::string> info;
};

inline State& state() {
  static State s;
  return s;
}

struct RequireFailed {};
struct Skipped {
  std::string why;
};

inline void report(bool ok, const char* macro, const char* expr, const char* file, int line) {
  ++state().assertions;
  if (ok) return;
  ++state().failures;
  std::fprintf(stderr, "%s:%d: FAILED: %s( %s )\n", file, line, macro, expr);
  for (const std::string& m : state().info) std::fprintf(stderr, "  with message: %s\n", m.c_str());
}

template <class F>
std::string to_message(F write) {
  std::ostringstream os;
  write(os);
  return os.str();
}

struct InfoScope {
  explicit InfoScope(std::string m) { state().info.push_back(std::move(m)); }
  ~InfoScope() { state().info.pop_back(); }
};

}  // namespace catch_min

#define CATCH_MIN_CAT2(a, b) a##b
#define CATCH_MIN_CAT(a, b) CATCH_MIN_CAT2(a, b)
#define CATCH_MIN_UNIQUE(base) CATCH_MIN_CAT(base, __LINE__)

#define CATCH_MIN_TEST_CASE2(fn, name, ...)                                               \
  static void fn();                                                                       \
  static const ::catch_min::Registrar CATCH_MIN_CAT(fn, _reg)(name, "" __VA_ARGS__, &fn); \
  static void fn()
#define TEST_CASE(...) CATCH_MIN_TEST_CASE2(CATCH_MIN_UNIQUE(catch_min_test_), __VA_ARGS__)

#define CHECK(...) ::catch_min::report(static_cast<bool>(__VA_ARGS__), "CHECK", #__VA_ARGS__, __FILE__, __LINE__)
#define CHECK_FALSE(...) \
  ::catch_min::report(!static_cast<bool>(__VA_ARGS__), "CHECK_FALSE", #__VA_ARGS__, __FILE__, __LINE__)
#define REQUIRE(...)                                                                          \
  do {                                                                                        \
    const bool catch_min_ok = static_cast<bool>(__VA_ARGS__);                                 \
    ::catch_min::report(catch_min_ok, "REQUIRE", #__VA_ARGS__, __FILE__, __LINE__);           \
    if (!catch_min_ok) throw ::catch_min::RequireFailed{};                                    \
  } while (0)
#define REQUIRE_FALSE(...) REQUIRE(!static_cast<bool>(__VA_ARGS__))

#define CATCH_MIN_THROWS_AS(macro, fatal, expr, type)                                     \
  do {                                                                                    \
    bool catch_min_ok = false;                                                            \
    try {                                                                                 \
      static_cast<void>(expr);                                                            \
    } catch (const type&) {                                                               \
      catch_min_ok = true;                                                                \
    } catch (...) {                                                                       \
    }                                                                                     \
    ::catch_min::report(catch_min_ok, macro, #expr ", " #type, __FILE__, __LINE__);       \
    if (fatal && !catch_min_ok) throw ::catch_min::RequireFailed{};                       \
  } while (0)
#define CHECK_THROWS_AS(expr, type) CATCH_MIN_THROWS_AS("CHECK_THROWS_AS", false, expr, type)
#define REQUIRE_THROWS_AS(expr, type) CATCH_MIN_THROWS_AS("REQUIRE_THROWS_AS", true, expr, type)
#define CHECK_NOTHROW(...)                                                              \
  do {                                                                                  \
    bool catch_min_ok = true;                                                           \
    try {                                                                               \
      static_cast<void>(__VA_ARGS__);                                                   \
    } catch (...) {                                                                     \
      catch_min_ok = false;                                                             \
    }                                                                                   \
    ::catch_min::report(catch_min_ok, "CHECK_NOTHROW", #__VA_ARGS__, __FILE__, __LINE__); \
  } while (0)

#define INFO(...)                                                 \
  const ::catch_min::InfoScope CATCH_MIN_UNIQUE(catch_min_info_)( \
      ::catch_min::to_message([&](std::ostream& catch_min_os) { catch_min_os << __VA_ARGS__; }))
#define SKIP(...) throw ::catch_min::Skipped{std::string("" __VA_ARGS__)}
#define SUCCEED(...) ::catch_min::report(true, "SUCCEED", "", __FILE__, __LINE__)
#define FAIL(...)                                                                 \
  do {                                                                            \
    ::catch_min::report(false, "FAIL", "" __VA_ARGS__, __FILE__, __LINE__);       \
    throw ::catch_min::RequireFailed{};                                           \
  } while (0)
