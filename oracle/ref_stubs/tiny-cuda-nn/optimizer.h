// Stub of tiny-cuda-nn's optimizer.h (oracle/_ref host build): nothing of it is used.
#pragma once
