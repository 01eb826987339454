// capi_adjoint.cpp — adjoint C-ABI (filled in with the adjoint pair).
#include "engine.h"
#include "runtime.h"
using namespace accel;
struct accel_adjoint { int dummy; };
extern "C" {
int accel_adjoint_create(accel_line*, int, int, int, const int32_t*, const int32_t*, const int32_t*, int, accel_adjoint**) { return fail(ACCEL_E_UNSUPPORTED, "adjoint not built"); }
int accel_adjoint_destroy(accel_adjoint*) { return ACCEL_OK; }
int accel_adjoint_forward(accel_adjoint*, const double*, double*) { return fail(ACCEL_E_UNSUPPORTED, "adjoint not built"); }
int accel_adjoint_backward(accel_adjoint*, const double*, double*, double*) { return fail(ACCEL_E_UNSUPPORTED, "adjoint not built"); }
}
