// Stub of tiny-cuda-nn's gpu_memory.h (oracle/_ref host build): nothing of it is used.
#pragma once
