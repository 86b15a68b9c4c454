/* Test infrastructure only: MATLAB's matrix.h is covered by the stand-in mex.h. */
#include "mex.h"
