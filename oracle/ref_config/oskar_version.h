/* Version macros for the reference library compiled by oracle/Makefile
 * (target ref_lib). The reference's own build writes this header from a
 * template with its release number; this test-only build has none, so the
 * values below only mark where the library came from. */
#ifndef OSKAR_VERSION_H_
#define OSKAR_VERSION_H_
#define OSKAR_VERSION 0x000000
#define OSKAR_VERSION_STR "reference (oracle build)"
#endif
