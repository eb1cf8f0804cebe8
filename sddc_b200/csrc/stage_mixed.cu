// Mixed form of the stage kernel: FP32 interpolation, fluxes and
// derivatives; FP64 state, RK update, pressure recovery and reductions.
#define SDDC_R float
#define SDDC_EXACT_FORM false
#define SDDC_LAUNCH launch_stage_mixed
#define SDDC_TRACE launch_trace_mixed
#define SDDC_VISC launch_visc_mixed
#include "stage_launch.inc"
