// hermite4-titan.h -- TEST INFRASTRUCTURE ONLY: SRC/hermite4.h includes this
// under -DCUDA_TITAN; it declares the noise-injecting CPU Gravity.
#pragma once
#define NOISE_GRAVITY_ORDER 4
#include "noise_gravity.inl"
