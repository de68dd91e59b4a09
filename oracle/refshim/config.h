/* Oracle build shim (test infrastructure only): the autoconf config.h the
 * reference sources include. */
#ifndef GX_ORACLE_CONFIG_H
#define GX_ORACLE_CONFIG_H
#define VERSION "oracle"
#define PACKAGE "mpifxcorr"
#define PACKAGE_VERSION "oracle"
#define HAVE_INTTYPES_H 1
#define HAVE_STDINT_H 1
#endif
