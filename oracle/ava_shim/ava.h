// Forwarding header of the CPU AVA stand-in (oracle test infrastructure).
#pragma once
#include "ava_shim.hpp"
