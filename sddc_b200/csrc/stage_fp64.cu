// FP64 form of the stage kernel with FMA contraction and reciprocals.
#define SDDC_R double
#define SDDC_EXACT_FORM false
#define SDDC_LAUNCH launch_stage_fp64
#define SDDC_TRACE launch_trace_fp64
#define SDDC_VISC launch_visc_fp64
#include "stage_launch.inc"
