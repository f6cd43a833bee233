// Exact flavour of the step kernel: built with --fmad=false and IEEE
// division/square root, so every cell rounds like the reference build.
#define SEIS_NS exact
#include "fd_step_impl.cuh"
