// nest's sod2d example as a callable function -- TEST INFRASTRUCTURE ONLY.
// examples/sod2d/sod2d.cpp is compiled where it lies; main() is renamed.
// Running it writes sod2d_*.dat into the current directory.
#ifndef NDEBUG
#define NDEBUG 1
#endif
#define main nest_ref_sod2d_main
#include "sod2d/sod2d.cpp"
#undef main

extern "C" int ref_sod2d_main(void) { return nest_ref_sod2d_main(); }
