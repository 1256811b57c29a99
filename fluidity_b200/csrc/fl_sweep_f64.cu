// FP64 instantiation of the sweep kernel.
#define FL_T double
#define FL_LAUNCH launch_sweep_f64
#define FL_TLOOP loop_transposes_f64
#include "fl_sweep_dispatch.inc"
