/* a_iso_3d_gpu -- drop-in for the reference a_iso_3d program
 * (a_iso_3d/a_iso_3d.c:224-804) running its time loop on the GPU.  Same
 * arguments and files; an extra "-P fp32|fp64|bfp16|fp16|bf16" picks the storage
 * precision. */
#include "../../include/seismod_gpu.h"

int main(int argc, char **argv) { return sm_a_iso_3d_main(argc, argv); }
