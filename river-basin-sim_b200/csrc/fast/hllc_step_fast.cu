// hllc_step_fast.cu -- the HLLC stage kernels of hllc_step.cu built a second time
// with fast arithmetic (RB_FAST_MATH: contracted multiply-adds, approximate
// division and square root), in namespace rb::fast. rb_set_arith_mode selects it.
#include "../hllc_step.cu"
