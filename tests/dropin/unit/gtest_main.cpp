// gtest_main.cpp -- runner for the tests registered through
// tests/dropin/unit/gtest/gtest.h: --gtest_filter=POS[-NEG] with ':'-separated
// '*' patterns on "Suite.Name", as GoogleTest's.  Test infrastructure only.
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "gtest/gtest.h"

namespace {

bool glob(const char* p, const char* s) {
  if (*p == '\0') return *s == '\0';
  if (*p == '*') return glob(p + 1, s) || (*s != '\0' && glob(p, s + 1));
  return *s != '\0' && (*p == '?' || *p == *s) && glob(p + 1, s + 1);
}

bool any_glob(const std::string& patterns, const std::string& name) {
  size_t a = 0;
  while (a <= patterns.size()) {
    size_t b = patterns.find(':', a);
    if (b == std::string::npos) b = patterns.size();
    if (glob(patterns.substr(a, b - a).c_str(), name.c_str())) return true;
    a = b + 1;
  }
  return false;
}

}  // namespace

int main(int argc, char** argv) {
  std::string pos = "*", neg;
  for (int i = 1; i < argc; ++i) {
    const char* kFlag = "--gtest_filter=";
    if (std::strncmp(argv[i], kFlag, std::strlen(kFlag)) == 0) {
      const std::string f = argv[i] + std::strlen(kFlag);
      const size_t dash = f.find('-');
      pos = dash == std::string::npos ? f : f.substr(0, dash);
      neg = dash == std::string::npos ? "" : f.substr(dash + 1);
      if (pos.empty()) pos = "*";
    }
  }
  int run = 0, failed = 0, skipped = 0;
  std::vector<std::string> failures;
  for (const auto& t : gtest_shim::registry()) {
    const std::string name = t.suite + "." + t.name;
    if (!any_glob(pos, name) || (!neg.empty() && any_glob(neg, name))) continue;
    ++run;
    gtest_shim::state() = gtest_shim::State{};
    std::printf("[ RUN      ] %s\n", name.c_str());
    std::fflush(stdout);
    try {
      t.fn();
    } catch (const std::exception& e) {
      gtest_shim::state().failed = true;
      std::printf("exception thrown from the test body: %s\n", e.what());
    } catch (...) {
      gtest_shim::state().failed = true;
      std::printf("unknown exception thrown from the test body\n");
    }
    if (gtest_shim::state().failed) {
      ++failed;
      failures.push_back(name);
      std::printf("[  FAILED  ] %s\n", name.c_str());
    } else if (gtest_shim::state().skipped) {
      ++skipped;
      std::printf("[  SKIPPED ] %s\n", name.c_str());
    } else {
      std::printf("[       OK ] %s\n", name.c_str());
    }
    std::fflush(stdout);
  }
  std::printf("[==========] %d tests ran: %d passed, %d failed, %d skipped.\n", run,
              run - failed - skipped, failed, skipped);
  for (const auto& f : failures) std::printf("[  FAILED  ] %s\n", f.c_str());
  return failed ? 1 : 0;
}
