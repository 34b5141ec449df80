// hermite8-titan.h -- TEST INFRASTRUCTURE ONLY: SRC/hermite8.h includes this
// under -DCUDA_TITAN; it declares the noise-injecting CPU Gravity.
#pragma once
#define NOISE_GRAVITY_ORDER 8
#include "noise_gravity.inl"
