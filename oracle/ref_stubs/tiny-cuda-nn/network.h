// Stub of tiny-cuda-nn's network.h (oracle/_ref host build): nothing of it is used.
#pragma once
