/* Shim config.h for compiling the reference's own sources in oracle/_ref. */
#ifndef BBT_SHIM_CONFIG_H
#define BBT_SHIM_CONFIG_H
#define PACKAGE_NAME "BIOBLOOMTOOLS"
#define PACKAGE_VERSION "2.3.4"
#define GIT_REVISION "2.3.4-oracle-shim"
#endif
