/* Global Arrays type-declaration header stand-in: nothing on the level-set
 * path uses its contents. */
#ifndef DCELL_ORACLE_MACDECLS_SHIM_H
#define DCELL_ORACLE_MACDECLS_SHIM_H
#endif
