// Stub of tiny-cuda-nn's encoding.h (oracle/_ref host build): nothing of it is used.
#pragma once
