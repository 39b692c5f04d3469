// Test infrastructure only: command-line front end of the CPU oracle, flag-compatible with the
// reference's dg_hdg_2d executable (dg_hdg_2d/src/main.cpp) plus --threads N.
#include "dgh_oracle.hpp"

int main(int argc, char **argv) { return oracle::run_main(argc, argv); }
