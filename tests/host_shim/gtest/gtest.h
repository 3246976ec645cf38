// Minimal stand-in for the googletest macros a Matter test file uses (TEST,
// ASSERT_NEAR, EXPECT_TRUE), so such a file builds against the B200 host
// Simulation without googletest.  Test infrastructure only.
//
// main() runs every registered test, or those named by --gtest_filter=A.B
// (exact names, ':'-separated), prints one "[ PASSED ]"/"[ FAILED ]" line per
// test and returns the number of failures.
#ifndef MATTER_GTEST_SHIM_H
#define MATTER_GTEST_SHIM_H

#include <cmath>
#include <cstring>
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace gtest_shim {

struct Case {
  std::string name;
  void (*fn)();
};

inline std::vector<Case>& registry() {
  static std::vector<Case> r;
  return r;
}

struct Failure {};

inline bool& current_failed() {
  static bool f = false;
  return f;
}

inline int add(const char* suite, const char* name, void (*fn)()) {
  registry().push_back({std::string(suite) + "." + name, fn});
  return 0;
}

inline void report(const char* file, int line, const std::string& what) {
  std::cout << file << ":" << line << ": Failure\n" << what << std::endl;
  current_failed() = true;
}

}  // namespace gtest_shim

#define TEST(suite, name)                                                                 \
  static void gtest_shim_##suite##_##name();                                              \
  static int gtest_shim_reg_##suite##_##name =                                            \
      gtest_shim::add(#suite, #name, &gtest_shim_##suite##_##name);                       \
  static void gtest_shim_##suite##_##name()

#define GTEST_SHIM_NEAR(a, b, tol, fatal)                                                 \
  do {                                                                                    \
    const double gs_a = (a), gs_b = (b), gs_t = (tol);                                    \
    if (!(std::fabs(gs_a - gs_b) <= gs_t)) {                                              \
      std::ostringstream gs_o;                                                            \
      gs_o.precision(17);                                                                 \
      gs_o << "|" #a " - " #b "| = " << std::fabs(gs_a - gs_b) << " > " << gs_t             \
           << " (" #a " = " << gs_a << ", " #b " = " << gs_b << ")";                      \
      gtest_shim::report(__FILE__, __LINE__, gs_o.str());                                 \
      if (fatal) throw gtest_shim::Failure();                                             \
    }                                                                                     \
  } while (0)

#define ASSERT_NEAR(a, b, tol) GTEST_SHIM_NEAR(a, b, tol, true)
#define EXPECT_NEAR(a, b, tol) GTEST_SHIM_NEAR(a, b, tol, false)

#define GTEST_SHIM_TRUE(c, fatal)                                                         \
  do {                                                                                    \
    if (!(c)) {                                                                           \
      gtest_shim::report(__FILE__, __LINE__, "expected true: " #c);                       \
      if (fatal) throw gtest_shim::Failure();                                             \
    }                                                                                     \
  } while (0)

#define EXPECT_TRUE(c) GTEST_SHIM_TRUE(c, false)
#define ASSERT_TRUE(c) GTEST_SHIM_TRUE(c, true)

int main(int argc, char** argv) {
  std::vector<std::string> only;
  for (int i = 1; i < argc; ++i) {
    const char* k = "--gtest_filter=";
    if (std::strncmp(argv[i], k, std::strlen(k)) == 0) {
      std::string s = argv[i] + std::strlen(k);
      size_t p = 0;
      while (p <= s.size()) {
        size_t q = s.find(':', p);
        if (q == std::string::npos) q = s.size();
        if (q > p) only.push_back(s.substr(p, q - p));
        p = q + 1;
      }
    }
  }
  int failures = 0, ran = 0;
  for (const auto& c : gtest_shim::registry()) {
    if (!only.empty()) {
      bool hit = false;
      for (const auto& o : only) hit |= (o == c.name);
      if (!hit) continue;
    }
    ++ran;
    gtest_shim::current_failed() = false;
    std::cout << "[ RUN      ] " << c.name << std::endl;
    try {
      c.fn();
    } catch (const gtest_shim::Failure&) {
    }
    if (gtest_shim::current_failed()) {
      ++failures;
      std::cout << "[  FAILED  ] " << c.name << std::endl;
    } else {
      std::cout << "[       OK ] " << c.name << std::endl;
    }
  }
  std::cout << "[==========] " << ran << " tests ran, " << failures << " failed." << std::endl;
  return failures;
}

#endif
