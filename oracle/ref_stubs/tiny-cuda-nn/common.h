// Stub of tiny-cuda-nn's common.h (oracle/_ref host build): the precision type only.
#pragma once
#include <cstdint>
namespace tcnn {
using network_precision_t = float;
}  // namespace tcnn
