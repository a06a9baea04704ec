// Stub (oracle/_ref host build): nothing of KiRaRay's window.h is used.
#pragma once
