// nest's sod1d example as a callable function -- TEST INFRASTRUCTURE ONLY.
// examples/sod1d/sod1d.cpp is compiled where it lies; main() is renamed.
// Running it writes sod_*.dat into the current directory.
#ifndef NDEBUG
#define NDEBUG 1
#endif
#define main nest_ref_sod1d_main
#include "sod1d/sod1d.cpp"
#undef main

extern "C" int ref_sod1d_main(void) { return nest_ref_sod1d_main(); }
