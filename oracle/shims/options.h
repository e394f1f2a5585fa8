/* Compile-only stand-in (oracle/_ref build only): included by optical_flow.h, unused. */
