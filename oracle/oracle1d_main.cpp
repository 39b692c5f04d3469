// Test infrastructure only: CLI of the 1D CPU oracle, flag-compatible with the reference's
// dg_hdg_1d program (dg_hdg_1d/src/config.cpp, main.cpp).
#include "dgh1d_oracle.hpp"
int main(int argc, char **argv) { return oracle1d::run_main(argc, argv); }
