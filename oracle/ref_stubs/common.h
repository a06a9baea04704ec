// Stub of KiRaRay's common.h for compiling reference helper functions on the host (test
// infrastructure for oracle/_ref). Declares only the macros the compiled reference code uses.
#pragma once
#include <cmath>
#include <cstdint>
#include <memory>
#define NAMESPACE_BEGIN(name) namespace name {
#define NAMESPACE_END(name) }
#define KRR_DEVICE_FUNCTION inline
#define KRR_CALLABLE inline
namespace nlohmann {
struct json {};
}  // namespace nlohmann
