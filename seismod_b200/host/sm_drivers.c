/* placeholder, replaced below */
#include "sm_host.h"
int sm_e_iso_main(int argc, char **argv) { (void)argc; (void)argv; return 1; }
int sm_a_iso_3d_main(int argc, char **argv) { (void)argc; (void)argv; return 1; }
