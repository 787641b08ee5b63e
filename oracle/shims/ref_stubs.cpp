// Stubs for two image-format writers/readers the reference dispatches to
// (bsoft/src/rwimg/rwimg.cpp:182, :390) whose sources need libjpeg / libtiff,
// neither of which is part of the reconstruction path or installed here.
#include "Bimage.h"
int writeJPEG(Bimage*, int) { return -1; }
int readEER(Bimage*, int, int, int) { return -1; }
