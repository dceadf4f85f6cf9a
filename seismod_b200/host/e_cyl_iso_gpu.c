/* e_cyl_iso_gpu -- drop-in for the reference e_cyl_iso program
 * (e_cyl_iso.c:277-885) running its time loop on the GPU.  Same arguments
 * and files; "-P fp32|fp64" picks the storage precision. */
#include "../../include/seismod_gpu.h"

int main(int argc, char **argv) { return sm_e_cyl_iso_main(argc, argv); }
