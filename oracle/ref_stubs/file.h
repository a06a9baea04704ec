// Stub (oracle/_ref host build): nothing of KiRaRay's file.h is used.
#pragma once
