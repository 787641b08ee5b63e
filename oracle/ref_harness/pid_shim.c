// A fixed process id for the reference programs.  breconstruct -mode 2 seeds
// random() with srandom(getpid()) (random_seed, bsoft/src/util/
// random_numbers.cpp:41-48); linked into a copy of breconstruct with
// -Wl,--wrap=getpid, this makes the seed the value of BSG_REF_PID, so that
// its random symmetric views are reproducible.  Test infrastructure only.
#include <stdlib.h>
#include <sys/types.h>

pid_t __real_getpid(void);

pid_t __wrap_getpid(void) {
    const char* s = getenv("BSG_REF_PID");
    return s ? (pid_t)atol(s) : __real_getpid();
}
