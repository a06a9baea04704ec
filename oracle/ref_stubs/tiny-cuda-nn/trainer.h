// Stub of tiny-cuda-nn's trainer.h (oracle/_ref host build): Trainer with its nested
// ForwardContext name, which the reference's type aliases refer to.
#pragma once
namespace tcnn {
template <typename T, typename PARAMS_T, typename COMPUTE_T>
class Trainer {
public:
    struct ForwardContext {};
};
}  // namespace tcnn
