// Fast flavour of the step kernel: the same source built with multiply-add
// contraction and approximate division (denormals kept), and the absorbing
// formulas' divisions by grid constants taken as products with reciprocals.
#define SEIS_NS fast
#define SEIS_FAST_MATH 1
#include "fd_step_impl.cuh"
