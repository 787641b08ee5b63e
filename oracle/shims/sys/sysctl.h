/* Empty stand-in for <sys/sysctl.h>, which glibc no longer ships.  The
 * reference includes it unconditionally (bsoft/src/util/utilities.cpp:10) but
 * only uses it behind a CTL_HW guard that is false on Linux. */
