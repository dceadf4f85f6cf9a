/*
 * The globals that the reference io_utils.c declares extern (io_utils.c:56-60)
 * and that each reference driver normally defines (e_iso.c:141-288).  Needed
 * only when the reference's own propagate.c / pml.c / src.c / io_utils.c are
 * linked into oracle/_ref/libref_eiso.so without a driver main().
 * Test infrastructure.
 */
int verbose = 0;
char *parFormat = "";
char *modelFormat = "";
char *srcFormat = "";
char *rcvFormat = "";
