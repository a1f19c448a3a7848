/* Global Arrays stand-in for compiling the reference's level-set path.
 * The oracle never fetches velocity through GA: callers fill the velocity
 * Grid directly, so these calls are link stubs that report failure. */
#ifndef DCELL_ORACLE_GA_SHIM_H
#define DCELL_ORACLE_GA_SHIM_H
void NGA_Get(int g_a, int lo[], int hi[], void *buf, int ld[]);
void NGA_Inquire(int g_a, int *type, int *ndim, int dims[]);
#endif
