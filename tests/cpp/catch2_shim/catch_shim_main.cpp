// The test runner of the Catch2 stand-in (main() of catch_test_macros.hpp).
#define CATCH_SHIM_MAIN
#include <catch2/catch_test_macros.hpp>
