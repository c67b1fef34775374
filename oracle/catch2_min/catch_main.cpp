// catch_main.cpp - runs the test cases registered through
// catch2/catch_test_macros.hpp (this directory). Test infrastructure.
//
//   <binary> [substring ...]   run the test cases whose name contains any of the
//                              substrings (all when none is given)
//
// Prints one line per test case (passed / FAILED / skipped) and a summary line
//   test cases: N | P passed | F failed | S skipped | A assertions
// and exits 0 when no test case failed, 1 otherwise.
#include <cstdio>
#include <cstring>
#include <exception>

#include "catch2/catch_test_macros.hpp"

int main(int argc, char** argv) {
  int n = 0, passed = 0, failed = 0, skipped = 0;
  for (const catch_min::TestCase& tc : catch_min::registry()) {
    bool selected = argc < 2;
    for (int i = 1; i < argc; ++i) selected = selected || std::strstr(tc.name, argv[i]) != nullptr;
    if (!selected) continue;
    ++n;
    catch_min::state().failures = 0;
    const char* verdict = "passed";
    std::string why;
    try {
      tc.fn();
    } catch (const catch_min::RequireFailed&) {
    } catch (const catch_min::Skipped& s) {
      verdict = "skipped";
      why = s.why;
    } catch (const std::exception& e) {
      ++catch_min::state().failures;
      std::fprintf(stderr, "%s: unexpected exception: %s\n", tc.name, e.what());
    } catch (...) {
      ++catch_min::state().failures;
      std::fprintf(stderr, "%s: unexpected exception\n", tc.name);
    }
    if (catch_min::state().failures > 0) verdict = "FAILED";
    if (std::strcmp(verdict, "passed") == 0) ++passed;
    else if (std::strcmp(verdict, "skipped") == 0) ++skipped;
    else ++failed;
    std::printf("[%s] %s%s%s\n", verdict, tc.name, why.empty() ? "" : ": ", why.c_str());
    std::fflush(stdout);
  }
  std::printf("test cases: %d | %d passed | %d failed | %d skipped | %ld assertions\n", n, passed,
              failed, skipped, catch_min::state().assertions);
  return failed == 0 ? 0 : 1;
}
