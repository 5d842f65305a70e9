/* Test-infrastructure shim: empty stand-in for CLAPACK's blaswrap.h. */
