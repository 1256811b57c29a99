// FP32 instantiation of the sweep kernel.
#define FL_T float
#define FL_LAUNCH launch_sweep_f32
#define FL_TLOOP loop_transposes_f32
#include "fl_sweep_dispatch.inc"
