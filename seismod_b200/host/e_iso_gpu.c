/* e_iso_gpu -- drop-in for the reference e_iso program (e_iso.c:290-699)
 * running its time loop on the GPU.  Same arguments and files; an extra
 * "-P fp32|fp64|bfp16|fp16|bf16" picks the storage precision. */
#include "../../include/seismod_gpu.h"

int main(int argc, char **argv) { return sm_e_iso_main(argc, argv); }
