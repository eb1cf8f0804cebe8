// FP64 exact form of the stage kernel: the reference's operations in its
// order, compiled with -fmad=false (no FMA contraction).
#define SDDC_R double
#define SDDC_EXACT_FORM true
#define SDDC_LAUNCH launch_stage_exact
#define SDDC_TRACE launch_trace_exact
#define SDDC_VISC launch_visc_exact
#include "stage_launch.inc"
