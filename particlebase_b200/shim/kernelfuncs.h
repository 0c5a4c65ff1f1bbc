// Drivers include kernelfuncs.h for the scalar type; the kernels themselves
// live in libparticlebase_b200.so.
#pragma once
#include "pb_shim.hh"
