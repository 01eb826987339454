// adjoint_params.h — parameter kinds of the adjoint, shared by host and device code.
#pragma once
#include <cstdint>

namespace accel {
namespace adj {
constexpr int kMaxParamsPerElem = 4;
enum ParamKind : int32_t { PK_B = 0, PK_A = 1, PK_QUADK = 2 };
}  // namespace adj
}  // namespace accel
