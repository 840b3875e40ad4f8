// catch2/catch_test_macros.hpp -- a small stand-in for the parts of Catch2
// v3.8.1 (pinned by the reference's CMakeLists.txt, absent from this image)
// that the reference's tests use: TEST_CASE, flat SECTIONs, REQUIRE,
// REQUIRE_FALSE, REQUIRE_NOTHROW, REQUIRE_THROWS_AS and REQUIRE_THAT.  It
// lets tests/*.cu|cpp of the reference compile unmodified against the
// drop-in headers.  Semantics kept from Catch2: a failed REQUIRE ends the
// current run of the test case; a test case with N sections runs N times,
// the k-th run entering only the k-th section.  One translation unit
// defines CATCH_SHIM_MAIN before including this header to get main().
#pragma once

#include <cstdio>
#include <cstring>
#include <exception>
#include <sstream>
#include <string>
#include <vector>

namespace catch_shim {

struct Failure {
  std::string what;
};

struct Case {
  const char* name;
  const char* tags;
  void (*fn)();
};

inline std::vector<Case>& registry() {
  static std::vector<Case> cases;
  return cases;
}

struct Registrar {
  Registrar(const char* name, const char* tags, void (*fn)()) {
    registry().push_back({name, tags, fn});
  }
};

struct Sections {
  int target = 0;  // the section this run enters
  int seen = 0;    // sections met so far in this run
};

inline Sections& sections() {
  static Sections s;
  return s;
}

inline bool enter_section() {
  Sections& s = sections();
  return s.seen++ == s.target;
}

[[noreturn]] inline void fail(const char* file, int line, const std::string& what) {
  std::ostringstream o;
  o << file << ":" << line << ": " << what;
  throw Failure{o.str()};
}

}  // namespace catch_shim

#define CATCH_SHIM_CAT2(a, b) a##b
#define CATCH_SHIM_CAT(a, b) CATCH_SHIM_CAT2(a, b)

#define TEST_CASE(name, tags)                                                        \
  static void CATCH_SHIM_CAT(catch_shim_case_, __LINE__)();                          \
  static catch_shim::Registrar CATCH_SHIM_CAT(catch_shim_reg_, __LINE__)(            \
      name, tags, &CATCH_SHIM_CAT(catch_shim_case_, __LINE__));                      \
  static void CATCH_SHIM_CAT(catch_shim_case_, __LINE__)()

#define SECTION(name) if (catch_shim::enter_section())

#define REQUIRE(...)                                                                 \
  do {                                                                               \
    if (!(__VA_ARGS__)) catch_shim::fail(__FILE__, __LINE__, "REQUIRE(" #__VA_ARGS__ ")"); \
  } while (0)

#define REQUIRE_FALSE(...)                                                           \
  do {                                                                               \
    if (__VA_ARGS__)                                                                 \
      catch_shim::fail(__FILE__, __LINE__, "REQUIRE_FALSE(" #__VA_ARGS__ ")");       \
  } while (0)

#define REQUIRE_NOTHROW(...)                                                         \
  do {                                                                               \
    try {                                                                            \
      __VA_ARGS__;                                                                   \
    } catch (const std::exception& catch_shim_e) {                                   \
      catch_shim::fail(__FILE__, __LINE__,                                           \
                       std::string("REQUIRE_NOTHROW(" #__VA_ARGS__ ") threw: ") +    \
                           catch_shim_e.what());                                     \
    } catch (...) {                                                                  \
      catch_shim::fail(__FILE__, __LINE__, "REQUIRE_NOTHROW(" #__VA_ARGS__ ") threw"); \
    }                                                                                \
  } while (0)

#define REQUIRE_THROWS_AS(expr, type)                                                \
  do {                                                                               \
    bool catch_shim_threw = false;                                                   \
    try {                                                                            \
      expr;                                                                          \
    } catch (const type&) {                                                          \
      catch_shim_threw = true;                                                       \
    } catch (...) {                                                                  \
      catch_shim::fail(__FILE__, __LINE__,                                           \
                       "REQUIRE_THROWS_AS(" #expr ", " #type ") threw another type"); \
    }                                                                                \
    if (!catch_shim_threw)                                                           \
      catch_shim::fail(__FILE__, __LINE__,                                           \
                       "REQUIRE_THROWS_AS(" #expr ", " #type ") did not throw");     \
  } while (0)

#define REQUIRE_THAT(arg, matcher)                                                   \
  do {                                                                               \
    const auto catch_shim_v = (arg);                                                 \
    const auto catch_shim_m = (matcher);                                             \
    if (!catch_shim_m.match(catch_shim_v)) {                                         \
      std::ostringstream catch_shim_o;                                               \
      catch_shim_o.precision(9);                                                     \
      catch_shim_o << "REQUIRE_THAT(" #arg ", " #matcher "): " << catch_shim_v << " "  \
                   << catch_shim_m.describe();                                       \
      catch_shim::fail(__FILE__, __LINE__, catch_shim_o.str());                      \
    }                                                                                \
  } while (0)

#ifdef CATCH_SHIM_MAIN
// Runs every registered test case (or those whose name contains argv[1]);
// one line per case: "PASS\t<name>" or "FAIL\t<name>\t<message>".  Exit
// status 1 when any case failed.
int main(int argc, char** argv) {
  const char* filter = argc > 1 ? argv[1] : nullptr;
  int passed = 0, failed = 0;
  for (const catch_shim::Case& c : catch_shim::registry()) {
    if (filter && !std::strstr(c.name, filter)) continue;
    std::string first_failure;
    for (int target = 0;; ++target) {
      catch_shim::sections() = catch_shim::Sections{target, 0};
      try {
        c.fn();
      } catch (const catch_shim::Failure& f) {
        if (first_failure.empty()) first_failure = f.what;
      } catch (const std::exception& e) {
        if (first_failure.empty()) first_failure = std::string("unexpected exception: ") + e.what();
      } catch (...) {
        if (first_failure.empty()) first_failure = "unexpected exception";
      }
      if (target + 1 >= catch_shim::sections().seen) break;
    }
    if (first_failure.empty()) {
      ++passed;
      std::printf("PASS\t%s\n", c.name);
    } else {
      ++failed;
      std::printf("FAIL\t%s\t%s\n", c.name, first_failure.c_str());
    }
    std::fflush(stdout);
  }
  std::printf("SUMMARY\t%d passed\t%d failed\n", passed, failed);
  return failed ? 1 : 0;
}
#endif
