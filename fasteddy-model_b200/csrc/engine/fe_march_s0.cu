// fe_march_s0.cu -- the i-marching stage kernel of RK stage 1 (both modes, every flavour).
#include "fasteddy_b200.h"
#include "fe_march_impl.cuh"

FE_MARCH_INSTANTIATE(0)
