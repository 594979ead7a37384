// li_step_fast.cu -- the local-inertial step kernels of li_step.cu built a second
// time with fast arithmetic (RB_FAST_MATH: contracted multiply-adds, approximate
// division and square root, __powf), in namespace rb::fast. rb_set_arith_mode
// selects it.
#include "../li_step.cu"
