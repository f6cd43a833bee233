// Fast flavour of the step kernel: the same source built with multiply-add
// contraction and approximate division (denormals kept).
#define SEIS_NS fast
#include "fd_step_impl.cuh"
