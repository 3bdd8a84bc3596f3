/* Build-time identity for the reference CLI compiled as a test oracle.
 * Prototype-only stand-in for the autotools-generated config.h. */
#ifndef OA_REF_CONFIG_H
#define OA_REF_CONFIG_H
#define PACKAGE_NAME "omicabelnomm"
#define PACKAGE_VERSION "reference-oracle"
#endif
