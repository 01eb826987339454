// kern_adjoint.cu — reverse-mode kernels (filled in with the adjoint pair).
#include "kernels.h"
