// Entry point of the conformance binary: runs every test registered through
// the minimal gtest header.
#include "gtest/gtest.h"

int main() { return ::gtm::run_all(); }
