// Stub of tiny-cuda-nn's cuda_graph.h (oracle/_ref host build): nothing of it is used.
#pragma once
