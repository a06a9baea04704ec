// Stub of tiny-cuda-nn's gpu_matrix.h (oracle/_ref host build): declarations only.
#pragma once
namespace tcnn {
template <typename T> class GPUMatrix;
}  // namespace tcnn
