// Opaque C-ABI handles shared by the ABI translation units.
#pragma once

#include "world.cuh"

struct PeWcsph {
    pe::World* world;
};
