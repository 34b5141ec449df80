// hermite6-titan.h -- TEST INFRASTRUCTURE ONLY: SRC/hermite6.h includes this
// under -DCUDA_TITAN; it declares the noise-injecting CPU Gravity.
#pragma once
#define NOISE_GRAVITY_ORDER 6
#include "noise_gravity.inl"
