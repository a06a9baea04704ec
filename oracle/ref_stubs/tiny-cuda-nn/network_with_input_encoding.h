// Stub of tiny-cuda-nn's network_with_input_encoding.h (oracle/_ref host build).
#pragma once
namespace tcnn {
template <typename T> class NetworkWithInputEncoding;
}  // namespace tcnn
